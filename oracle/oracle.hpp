// oracle.hpp — FP64 CPU restatement of EulerianFSI.jl's IMEX fractional step.
//
// TEST INFRASTRUCTURE ONLY.  This oracle is the checker the GPU path is compared
// against; nothing in the product path links or calls it.  It follows the
// reference Julia sources function by function (citations are file:line within
// the EulerianFSI.jl project) with 0-based indices: a Julia loop index k maps to
// k-1 here.  Arrays are column-major (x index fastest) like Julia matrices.
//
// Parity pinning: Julia is not available, so the oracle is pinned by the
// reference's own known-answer tests (test/runtests.jl, test/growth_tests.jl),
// restated in tests/test_oracle_known_answers.py.  Full-step outputs have no
// reference golden vectors; the linear solves are converged to ~1e-13 so the
// result is the unique solution of each discrete system.
#pragma once

#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../include/efsi.h"

namespace ora {

struct Err : std::runtime_error {
    int code;
    Err(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
[[noreturn]] inline void arg_error(const std::string& m) { throw Err(EFSI_ARG, m); }
[[noreturn]] inline void dim_error(const std::string& m) { throw Err(EFSI_DIM, m); }
[[noreturn]] inline void solve_error(const std::string& m) { throw Err(EFSI_SOLVE, m); }
[[noreturn]] inline void domain_error(const std::string& m) { throw Err(EFSI_DOMAIN, m); }

// Column-major 2-D field.
struct F2 {
    int nx = 0, ny = 0;
    std::vector<double> a;
    F2() = default;
    F2(int nx_, int ny_, double v = 0.0) : nx(nx_), ny(ny_), a((size_t)nx_ * ny_, v) {}
    double& operator()(int i, int j) { return a[(size_t)i + (size_t)j * nx]; }
    double operator()(int i, int j) const { return a[(size_t)i + (size_t)j * nx]; }
    size_t size() const { return a.size(); }
};

// MeshMetrics (MeshGeneration.jl:41-73).
struct Mesh {
    int Nx = 0, Ny = 0;
    double Lx = 0, Ly = 0;
    bool px = false, py = false;
    std::vector<double> dx_f, dx_c, dy_f, dy_c;
    std::vector<double> wL_c2fx, wR_c2fx, wB_c2fy, wT_c2fy;
    std::vector<double> wL_f2cx, wR_f2cx, wB_f2cy, wT_f2cy;
    std::vector<double> dxw, dxe, dys, dyn;  // dx_west/east_corner, dy_south/north_corner
};

// One side of a BoundaryConditionSetup (BoundaryConditions.jl:23-72).
struct Side {
    int type = EFSI_BC_NEUMANN;
    std::vector<double> value, neumann;
    std::vector<uint8_t> mask;
    double val(int k) const;             // boundary_value / mixed_dirichlet_value / backflow_value
    double neu(int k) const;             // mixed_neumann_value
    bool is_dir(int k) const;            // mixed_is_dirichlet
};
struct BCS {
    Side s[4];  // left, right, bottom, top
    const Side& left() const { return s[0]; }
    const Side& right() const { return s[1]; }
    const Side& bottom() const { return s[2]; }
    const Side& top() const { return s[3]; }
    bool periodic_x() const { return s[0].type == EFSI_BC_PERIODIC; }
    bool periodic_y() const { return s[2].type == EFSI_BC_PERIODIC; }
    bool has_dirichlet() const;
};

Mesh make_mesh(const efsi_mesh& m);
BCS make_bcs(const efsi_bc_setup& b, int n_lr, int n_bt, const char* name);

// ---- Operators.jl -----------------------------------------------------------
F2 interp_c2fx(const F2& f, const Mesh& m);                  // Operators.jl:110-133
F2 interp_c2fy(const F2& f, const Mesh& m);                  // Operators.jl:136-159
F2 interp_c2corners(const F2& f, const Mesh& m);             // Operators.jl:162-185
void scalar_gradient(const F2& f, const Mesh& m, const BCS& bc, F2& gx, F2& gy);  // :189-356, :395-404
F2 divergence(const F2& U, const F2& V, const Mesh& m);      // Operators.jl:407-425
void velocity_gradient(const F2& U, const F2& V, const Mesh& m, const BCS& bu, const BCS& bv,
                       F2& dudx, F2& dudy, F2& dvdx, F2& dvdy);               // :431-586
void symmetric_stress_divergence(const F2& Txx, const F2& Tyy, const F2& Txy, const Mesh& m,
                                 F2& Fx, F2& Fy);                              // :620-735
F2 diffusion_apply(const F2& c, const F2& D, const Mesh& m, const BCS& bc);   // :361-384 (+:1115)
void diffusion_matrix_apply(const F2& c, const F2& D, const Mesh& m, const BCS& bc, F2& out);
// Viscous affine operator (Operators.jl:848-1083) applied to a compact vector.
void viscous_apply(const std::vector<double>& x, const F2& mu, const Mesh& m, const BCS& bu,
                   const BCS& bv, bool with_boundary, std::vector<double>& out);
void velocity_dirichlet_data(const Mesh& m, const BCS& bu, const BCS& bv,
                             std::vector<int>& idx, std::vector<double>& val);  // :1085-1110

// ---- physics ----------------------------------------------------------------
struct Models;
void material_convection(const F2& U, const F2& V, const F2& S, const Mesh& m, const BCS& bu,
                         const BCS& bv, F2& Cu, F2& Cv);                        // MomentumTransport.jl:303-337
F2 phase_field_rhs(const efsi_models& md, const F2& U, const F2& V, const F2& phi, const F2& S,
                   const Mesh& m, const BCS& bphi);
F2 uwcdi_strang_step(const efsi_models& md, const F2& U, const F2& V, const F2& phi, double dt,
                     const Mesh& m, const BCS& bphi, bool x_first);             // PhaseFieldMethods.jl:810-850
void structure_tensor_rhs(const F2& sxx, const F2& syy, const F2& sxy, const F2& U, const F2& V,
                          const F2& Kxx, const F2& Kxy, const F2& Kyx, const F2& Kyy,
                          const efsi_models& md, const efsi_numerics& nu, const Mesh& m,
                          const BCS* bsig, const BCS& bu, const BCS& bv, const F2& phi,
                          F2& rxx, F2& ryy, F2& rxy);                           // StructureTensor.jl:377-463
void sigma_log_product_2d(double a, double d, double b, double& oxx, double& oyy, double& oxy);
void structure_extension_rhs(const efsi_numerics& nu, const F2& sxx, const F2& syy, const F2& sxy,
                             const F2& phi, F2& rxx, F2& ryy, F2& rxy);         // :469-551
int apply_structure_extension(const efsi_numerics& nu, F2& sxx, F2& syy, F2& sxy, const F2& phi);
struct SigmaDiag { double min_det, max_abs_det_err, min_eig; long long non_spd; };
SigmaDiag structure_tensor_diagnostics(const F2& sxx, const F2& syy, const F2& sxy);  // :627-662
void capillary_force(const efsi_models& md, const F2& phi, const Mesh& m, const BCS& bphi,
                     F2& Fx, F2& Fy);                                           // Capillarity.jl:123-188
void body_force(const efsi_models& md, double t, const Mesh& m, F2& Fx, F2& Fy);  // TransportConstitutive.jl:369-397
void viscosity_field(const efsi_models& md, const F2& phi, F2& out);           // :131-165
void diffusivity_field(const efsi_models& md, const F2& phi, F2& out);         // :217-240
void resource_sink(const efsi_models& md, const F2& phi, const F2& c, F2& out);  // :279-299
void growth_source(const efsi_models& md, const F2& phi, const F2& c, F2& G);  // GrowthModels.jl:214-250
void growth_tensor(const efsi_models& md, const F2& G, F2& Kxx, F2& Kxy, F2& Kyx, F2& Kyy);  // :268-318
double growth_trace_error(const F2& G, const F2& Kxx, const F2& Kyy);          // :336-352
F2 resource_explicit_rhs(const F2& U, const F2& V, const F2& c, const F2& sink, const Mesh& m,
                         const BCS& bc);                                        // ResourceTransport.jl:292-342
void relaxation_rhs(const efsi_models& md, double sxx, double syy, double sxy,
                    double& rxx, double& ryy, double& rxy);                    // StructuralConstitutive.jl:61-85

// ---- solvers ----------------------------------------------------------------
// Cavity-driver diagnostics (run_sugiyama_lid_driven_cavity.jl:484-828).
void state_diagnostics(const Mesh& m, const BCS& bphi, const F2& U, const F2& V, const F2& phi, const F2& sxx,
                       const F2& syy, const F2& sxy, const efsi_diag_config& cfg, efsi_diagnostics& out);
// tensor_cell_diagnostics_2d (BenchmarkUtilities.jl:62-87): det, det-1, lambda_min, lambda_max, stress.
void tensor_cell_diagnostics(double sxx, double syy, double sxy, double phi, double modulus, double out[5]);

struct Projector;
struct ProjOut { double linear_relative_residual, constraint_linf, constraint_l2, compatibility_defect; int iters; };
Projector* make_projector(const Mesh& m, const BCS& bq);
void free_projector(Projector* p);
ProjOut project(Projector* p, F2& U, F2& V, const F2& target, F2& correction, double reltol,
                int maxiter);                                                  // Projection.jl:170-307
// x <- solution of A x = b by restarted BiCGSTAB to relative residual tol.
template <class Op>
int bicgstab(const Op& A, const std::vector<double>& b, std::vector<double>& x, double tol, int maxiter);

}  // namespace ora
