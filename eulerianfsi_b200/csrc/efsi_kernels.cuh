// efsi_kernels.cuh — launch wrappers of the IMEX-step kernels (host side).
#pragma once

#include "efsi_common.cuh"

namespace efsi {

// Buffers of one stage state (device pointers).
struct StageFields {
    const double *U, *V, *phi, *c, *sxx, *syy, *sxy, *G;
};

// ---- efsi_ops.cu ----
void launch_prepare_step(const Params& P, const double* U, const double* V, const double* phi,
                         const double* c, const double* sxx, const double* syy, const double* sxy,
                         double* sxn, double* syn, double* sxyn, DevStatus* st, cudaStream_t s);
void launch_combine_scalars(const Params& P, int stage, const double* dt, const double* phin,
                            const double* sxn, const double* syn, const double* sxyn, const double* cn,
                            double* const* Ephi, double* const* Exx, double* const* Eyy,
                            double* const* Exy, double* const* Ec, double* const* Ic, double* phis,
                            double* sxs, double* sys, double* sxys, double* cs_or_rhs, cudaStream_t s);
void launch_velocity_rhs(const Params& P, int stage, const double* dt, const double* Un, const double* Vn,
                         double* const* Eu, double* const* Ev, double* const* Iu, double* const* Iv,
                         const double* phis, double* rhs_u, double* rhs_v, cudaStream_t s);
void launch_growth(const Params& P, const double* phi, const double* c, double* G, double* trace_max,
                   const RedSlot& rs, cudaStream_t s);
void launch_stage1_check(const Params& P, const double* U, const double* V, const double* G,
                         double* out_linf, const RedSlot& rs, DevStatus* st, cudaStream_t s);
void launch_momentum_rhs(const Params& P, double t, const StageFields& f, const double* kappa,
                         double* Eu, double* Ev, DevStatus* st, cudaStream_t s);
void launch_momentum_full(const Params& P, double t, const StageFields& f, const double* kappa,
                          double* Fx, double* Fy, DevStatus* st, cudaStream_t s);
void launch_capillary_curvature(const Params& P, const double* phi, double* smooth_a, double* smooth_b,
                                double* kappa, cudaStream_t s);
void launch_viscous_apply(const Params& P, const double* U, const double* V, const double* phi,
                          double* Iu, double* Iv, cudaStream_t s);
void launch_structure_rhs(const Params& P, const StageFields& f, double* Exx, double* Eyy, double* Exy,
                          DevStatus* st, cudaStream_t s);
void launch_resource_rhs(const Params& P, const StageFields& f, double* Ec, double* Ic, DevStatus* st,
                         cudaStream_t s);
void launch_finalize(const Params& P, const double* Us, const double* Vs, const double* phis,
                     const double* cs, const double* sxs, const double* sys, const double* sxys, double* U,
                     double* V, double* phi, double* c, double* sxx, double* syy, double* sxy,
                     double* report6, long long* nonspd, const RedSlot& rmin, const RedSlot& rmax,
                     const DevStatus* st, cudaStream_t s);
void launch_phase_rhs(const Params& P, const StageFields& f, const double* gamma_eff, double* Ephi,
                      DevStatus* st, cudaStream_t s);
// One directional sweep of uwcdi_strang_step (axis 1 = x, 2 = y), out = phi - h div(F).
void launch_strang_sweep(const Params& P, const double* U, const double* V, const double* phi, double* out, int axis,
                         double h, DevStatus* st, cudaStream_t s);
void launch_umax(const Params& P, const double* U, const double* V, double* out, const RedSlot& rs,
                 cudaStream_t s);
void launch_copy(double* dst, const double* src, size_t n, cudaStream_t s);

}  // namespace efsi
