// efsi_ops.cu — explicit kernels of the IMEX fractional step on sm_100a:
// step preparation, stage combination, growth fields, momentum forcing, the
// compact viscous operator, structure-tensor and resource tendencies, and the
// final commit with the StepReport reductions.
//
// All of these are HBM-bound stencils (well under 10 FP64 flop/byte); one thread
// owns one cell / MAC face and reads its neighbours through L1, so every field
// is streamed once per kernel in x-fastest, warp-coalesced rows.
#include <algorithm>
#include <cmath>

#include "efsi_device.cuh"
#include "efsi_kernels.cuh"

namespace efsi {

static constexpr int BX = 32, BY = 8;
static inline dim3 grid2(int nx, int ny) { return dim3((nx + BX - 1) / BX, (ny + BY - 1) / BY); }

// Tableaux (TimeIntegrationIMEX.jl:74-90).
__constant__ double c_AE[4][4] = {{0, 0, 0, 0}, {8.0 / 15, 0, 0, 0}, {1.0 / 4, 5.0 / 12, 0, 0}, {1.0 / 4, 0, 3.0 / 4, 0}};
__constant__ double c_AI[4][4] = {{0, 0, 0, 0}, {4.0 / 15, 4.0 / 15, 0, 0}, {4.0 / 15, 1.0 / 3, 1.0 / 15, 0},
                                  {4.0 / 15, 1.0 / 3, 7.0 / 30, 1.0 / 6}};

// ---- prepare: validation and time-n structure-tensor reset ---------------------------------
__device__ __forceinline__ bool ext_reset(const efsi_numerics& nu, double phi) {  // StructureTensor.jl:553-613
    if (nu.structure_extension == EFSI_EXT_IDENTITY_OUTSIDE) return phi < nu.extension_cutoff;
    if (nu.structure_extension == EFSI_EXT_GEOMETRIC) return nu.extension_cutoff > 0.0 && phi < nu.extension_cutoff;
    return false;
}

__global__ void k_prepare(Params P, const double* __restrict__ U, const double* __restrict__ V,
                          const double* __restrict__ phi, const double* __restrict__ c,
                          const double* __restrict__ sxx, const double* __restrict__ syy,
                          const double* __restrict__ sxy, double* sxn, double* syn, double* sxyn,
                          DevStatus* st) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    if (i <= Nx && j < Ny) {
        double u = U[uidx(i, j, Nx)];
        if (!isfinite(u)) raise_err(st, DE_NONFINITE_STATE, 0, i, j, u);
    }
    if (i < Nx && j <= Ny) {
        double v = V[vidx(i, j, Nx)];
        if (!isfinite(v)) raise_err(st, DE_NONFINITE_STATE, 1, i, j, v);
    }
    if (i < Nx && j < Ny) {
        size_t k = cidx(i, j, Nx);
        double p = phi[k], r = c[k], a = sxx[k], d = syy[k], b = sxy[k];
        if (!isfinite(p)) raise_err(st, DE_NONFINITE_STATE, 2, i, j, p);
        if (!isfinite(r)) raise_err(st, DE_NONFINITE_STATE, 3, i, j, r);
        if (!isfinite(a)) raise_err(st, DE_NONFINITE_STATE, 4, i, j, a);
        if (!isfinite(d)) raise_err(st, DE_NONFINITE_STATE, 5, i, j, d);
        if (!isfinite(b)) raise_err(st, DE_NONFINITE_STATE, 6, i, j, b);
        if (ext_reset(P.nu, p)) { a = 1.0; d = 1.0; b = 0.0; }
        sxn[k] = a; syn[k] = d; sxyn[k] = b;
    }
}

void launch_prepare_step(const Params& P, const double* U, const double* V, const double* phi, const double* c,
                         const double* sxx, const double* syy, const double* sxy, double* sxn, double* syn,
                         double* sxyn, DevStatus* st, cudaStream_t s) {
    k_prepare<<<grid2(P.g.Nx + 1, P.g.Ny + 1), dim3(BX, BY), 0, s>>>(P, U, V, phi, c, sxx, syy, sxy, sxn, syn,
                                                                     sxyn, st);
}

// ---- stage combination (TimeIntegrationIMEX.jl:716-774) ---------------------------------------
struct HistPtrs {
    const double* p[3];
};

__global__ void k_combine_scalars(Params P, int s, const double* __restrict__ dtp, const double* __restrict__ phin,
                                  const double* __restrict__ sxn, const double* __restrict__ syn,
                                  const double* __restrict__ sxyn, const double* __restrict__ cn, HistPtrs Ephi,
                                  HistPtrs Exx, HistPtrs Eyy, HistPtrs Exy, HistPtrs Ec, HistPtrs Ic, double* phis,
                                  double* sxs, double* sys, double* sxys, double* cs) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx;
    if (i >= Nx || j >= P.g.Ny) return;
    const double dt = *dtp;
    size_t k = cidx(i, j, Nx);
    double p = phin[k], a = sxn[k], d = syn[k], b = sxyn[k], r = cn[k];
    for (int q = 0; q < s; ++q) {
        double ae = c_AE[s][q];
        if (ae != 0.0) {
            double w = dt * ae;
            p += w * Ephi.p[q][k];
            a += w * Exx.p[q][k];
            d += w * Eyy.p[q][k];
            b += w * Exy.p[q][k];
        }
        double ai = c_AI[s][q];
        if (cs && (ae != 0.0 || ai != 0.0) && Ec.p[q])
            r += dt * (ae * Ec.p[q][k] + ai * (Ic.p[q] ? Ic.p[q][k] : 0.0));
    }
    if (ext_reset(P.nu, p)) { a = 1.0; d = 1.0; b = 0.0; }
    phis[k] = p; sxs[k] = a; sys[k] = d; sxys[k] = b;
    if (cs) {
        if (P.md.diffusivity != EFSI_DIFF_NONE) {
            // + alpha * boundary of the diffusion operator (:759); the boundary vector
            // is nonzero only in cells touching a Dirichlet / Neumann-data face.
            double alpha = dt * c_AI[s][s];
            const int Ny = P.g.Ny;
            double bnd = 0.0;
            double D = diffusivity(P.md, p);
            // x faces
            if (!P.g.px) {
                if (i == 0) {
                    const SideD& sd = P.bc.s[LEFT];
                    double g;
                    if (bdir(sd, j)) g = -bval(sd, j) / (0.5 * P.g.hx);
                    else if (sd.type == EFSI_BC_NEUMANN) g = -bval(sd, j);
                    else if (sd.type == EFSI_BC_MIXED) g = -bneu(sd, j);
                    else g = 0.0;
                    bnd += -(D * g) * P.g.ihx;
                }
                if (i == Nx - 1) {
                    const SideD& sd = P.bc.s[RIGHT];
                    double g;
                    if (bdir(sd, j)) g = bval(sd, j) / (0.5 * P.g.hx);
                    else if (sd.type == EFSI_BC_NEUMANN) g = bval(sd, j);
                    else if (sd.type == EFSI_BC_MIXED) g = bneu(sd, j);
                    else g = 0.0;
                    bnd += (D * g) * P.g.ihx;
                }
            }
            if (!P.g.py) {
                if (j == 0) {
                    const SideD& sd = P.bc.s[BOTTOM];
                    double g;
                    if (bdir(sd, i)) g = -bval(sd, i) / (0.5 * P.g.hy);
                    else if (sd.type == EFSI_BC_NEUMANN) g = -bval(sd, i);
                    else if (sd.type == EFSI_BC_MIXED) g = -bneu(sd, i);
                    else g = 0.0;
                    bnd += -(D * g) * P.g.ihy;
                }
                if (j == Ny - 1) {
                    const SideD& sd = P.bc.s[TOP];
                    double g;
                    if (bdir(sd, i)) g = bval(sd, i) / (0.5 * P.g.hy);
                    else if (sd.type == EFSI_BC_NEUMANN) g = bval(sd, i);
                    else if (sd.type == EFSI_BC_MIXED) g = bneu(sd, i);
                    else g = 0.0;
                    bnd += (D * g) * P.g.ihy;
                }
            }
            r += alpha * bnd;
        }
        cs[k] = r;
    }
}

void launch_combine_scalars(const Params& P, int stage, const double* dt, const double* phin, const double* sxn,
                            const double* syn, const double* sxyn, const double* cn, double* const* Ephi,
                            double* const* Exx, double* const* Eyy, double* const* Exy, double* const* Ec,
                            double* const* Ic, double* phis, double* sxs, double* sys, double* sxys,
                            double* cs_or_rhs, cudaStream_t s) {
    HistPtrs a{}, b{}, c{}, d{}, e{}, f{};
    for (int q = 0; q < 3; ++q) {
        a.p[q] = Ephi[q]; b.p[q] = Exx[q]; c.p[q] = Eyy[q]; d.p[q] = Exy[q];
        e.p[q] = Ec ? Ec[q] : nullptr; f.p[q] = Ic ? Ic[q] : nullptr;
    }
    k_combine_scalars<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, stage, dt, phin, sxn, syn, sxyn, cn, a, b, c,
                                                                   d, e, f, phis, sxs, sys, sxys, cs_or_rhs);
}

// Viscous boundary vector entries (Operators.jl:958-1080) at compact rows.
__device__ __forceinline__ void visc_boundary(const Params& P, const MuField& mu, int i, int j, double& bu,
                                              double& bv) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const double hx = P.g.hx, hy = P.g.hy;
    bu = 0.0; bv = 0.0;
    if (!P.g.px && i == Nx - 1) bu += (2.0 * mu.c(i, j) * (bval(P.bu.s[RIGHT], j) * P.g.ihx)) * P.g.ihx;
    if (!P.g.py && j == Ny - 1) bv += (2.0 * mu.c(i, j) * (bval(P.bv.s[TOP], i) * P.g.ihy)) * P.g.ihy;
    if (!P.g.py) {
        if (j == 0 && P.bu.s[BOTTOM].type == EFSI_BC_DIRICHLET)
            bu += mu.k(i, 0) / (hy * (0.5 * hy)) * bval(P.bu.s[BOTTOM], i);
        if (j == Ny - 1 && P.bu.s[TOP].type == EFSI_BC_DIRICHLET)
            bu += mu.k(i, Ny) / (hy * (0.5 * hy)) * bval(P.bu.s[TOP], i);
    }
    if (!P.g.px) {
        if (i == 0 && P.bv.s[LEFT].type == EFSI_BC_DIRICHLET)
            bv += mu.k(0, j) / (hx * (0.5 * hx)) * bval(P.bv.s[LEFT], j);
        if (i == Nx - 1 && P.bv.s[RIGHT].type == EFSI_BC_DIRICHLET)
            bv += mu.k(Nx, j) / (hx * (0.5 * hx)) * bval(P.bv.s[RIGHT], j);
    }
}

__global__ void k_velocity_rhs(Params P, int s, const double* __restrict__ dtp, const double* __restrict__ Un,
                               const double* __restrict__ Vn, HistPtrs Eu, HistPtrs Ev, HistPtrs Iu, HistPtrs Iv,
                               const double* __restrict__ phis, double* rhs_u, double* rhs_v) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    if (i >= Nx || j >= Ny) return;
    const double dt = *dtp;
    size_t k = cidx(i, j, Nx);
    double ru = Un[uidx(i, j, Nx)], rv = Vn[vidx(i, j, Nx)];
    for (int q = 0; q < s; ++q) {  // TimeIntegrationIMEX.jl:777-784
        double ae = c_AE[s][q], ai = c_AI[s][q];
        if (ae != 0.0 || ai != 0.0) {
            ru += dt * (ae * Eu.p[q][k] + ai * Iu.p[q][k]);
            rv += dt * (ae * Ev.p[q][k] + ai * Iv.p[q][k]);
        }
    }
    if (P.md.viscosity != EFSI_VISC_NONE) {  // :790-792
        MuField mu = make_mu(P, phis);
        double alpha = dt * c_AI[s][s];
        double bu, bv;
        visc_boundary(P, mu, i, j, bu, bv);
        ru += alpha * bu;
        rv += alpha * bv;
    }
    rhs_u[k] = ru;
    rhs_v[k] = rv;
}

void launch_velocity_rhs(const Params& P, int stage, const double* dt, const double* Un, const double* Vn,
                         double* const* Eu, double* const* Ev, double* const* Iu, double* const* Iv,
                         const double* phis, double* rhs_u, double* rhs_v, cudaStream_t s) {
    HistPtrs a{}, b{}, c{}, d{};
    for (int q = 0; q < 3; ++q) { a.p[q] = Eu[q]; b.p[q] = Ev[q]; c.p[q] = Iu[q]; d.p[q] = Iv[q]; }
    k_velocity_rhs<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, stage, dt, Un, Vn, a, b, c, d, phis, rhs_u,
                                                                rhs_v);
}

// ---- growth fields (TimeIntegrationIMEX.jl:842-865) ---------------------------------------------
__global__ void k_growth(Params P, const double* __restrict__ phi, const double* __restrict__ c, double* G,
                         double* trace_max, RedSlot rs) {
    __shared__ double sh[32];
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx;
    double te[1] = {0.0};
    if (i < Nx && j < P.g.Ny) {
        size_t k = cidx(i, j, Nx);
        double g = growth_G(P.md, phi[k], c[k]);
        G[k] = g;
        double kxx, kxy, kyx, kyy;
        growth_K(P.md, g, kxx, kxy, kyx, kyy);
        te[0] = fabs(kxx + kyy - g);
    }
    double tot[1];
    if (grid_reduce<1, true>(te, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0)
        *trace_max = fmax(*trace_max, tot[0]);
}

void launch_growth(const Params& P, const double* phi, const double* c, double* G, double* trace_max,
                   const RedSlot& rs, cudaStream_t s) {
    k_growth<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, phi, c, G, trace_max, rs);
}

// ---- stage-1 constraint (TimeIntegrationIMEX.jl:1111-1127) ------------------------------------
__global__ void k_stage1_check(Params P, const double* __restrict__ U, const double* __restrict__ V,
                               const double* __restrict__ G, double* out_linf, RedSlot rs, DevStatus* st) {
    __shared__ double sh[64];
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx;
    double v[2] = {0.0, 0.0};
    if (i < Nx && j < P.g.Ny) {
        double div = (U[uidx(i + 1, j, Nx)] - U[uidx(i, j, Nx)]) * P.g.ihx +
                     (V[vidx(i, j + 1, Nx)] - V[vidx(i, j, Nx)]) * P.g.ihy;
        double g = G ? G[cidx(i, j, Nx)] : 0.0;
        v[0] = fabs(div - g);
        v[1] = fabs(g);
    }
    double tot[2];
    if (grid_reduce<2, true>(v, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        *out_linf = fmax(*out_linf, tot[0]);
        if (P.nu.check_stage1_constraint) {
            double tol = P.nu.stage1_constraint_atol + P.nu.stage1_constraint_rtol * fmax(tot[1], 1.0);
            if (!(tot[0] <= tol)) raise_err(st, DE_STAGE1_CONSTRAINT, 1, -1, -1, tot[0]);
        }
    }
}

void launch_stage1_check(const Params& P, const double* U, const double* V, const double* G, double* out_linf,
                         const RedSlot& rs, DevStatus* st, cudaStream_t s) {
    k_stage1_check<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, U, V, G, out_linf, rs, st);
}

// ---- momentum forcing (TimeIntegrationIMEX.jl:959-985) --------------------------------------------
struct Cells {
    const double *phi, *sxx, *syy, *sxy, *G;
};

// Combined cell stress phi*tau_e + growth-viscous stress (TimeIntegrationIMEX.jl:903-942);
// both enter through the same linear symmetric_stress_divergence.
__device__ __forceinline__ void cell_stress(const Params& P, const Cells& f, int i, int j, double& txx,
                                            double& tyy, double& txy) {
    size_t k = cidx(i, j, P.g.Nx);
    txx = tyy = txy = 0.0;
    double phi = f.phi[k];
    if (P.md.elastic_stress == EFSI_ELASTIC_LINEAR) {
        double g = P.md.elastic_coefficient;
        txx = phi * (g * (f.sxx[k] - 1.0));
        tyy = phi * (g * (f.syy[k] - 1.0));
        txy = phi * (g * f.sxy[k]);
    }
    if (P.md.viscosity != EFSI_VISC_NONE && f.G) {
        double G = f.G[k], kxx, kxy, kyx, kyy;
        growth_K(P.md, G, kxx, kxy, kyx, kyy);
        double mu = viscosity(P.md, phi);
        txx += -2.0 * mu * kxx;
        tyy += -2.0 * mu * kyy;
        txy += -mu * (kxy + kyx);
    }
}
__device__ __forceinline__ double cell_txx(const Params& P, const Cells& f, int i, int j) {
    double a, b, c; cell_stress(P, f, i, j, a, b, c); return a;
}
__device__ __forceinline__ double cell_tyy(const Params& P, const Cells& f, int i, int j) {
    double a, b, c; cell_stress(P, f, i, j, a, b, c); return b;
}
__device__ __forceinline__ double cell_txy(const Params& P, const Cells& f, int i, int j) {
    double a, b, c; cell_stress(P, f, i, j, a, b, c); return c;
}

// Txy on x-face i at row r (Operators.jl:770-789, linear extrapolation at walls).
__device__ __forceinline__ double txy_xface(const Params& P, const Cells& f, int i, int r) {
    const int Nx = P.g.Nx;
    if (P.g.px) {
        if (i == 0 || i == Nx) return 0.5 * (cell_txy(P, f, Nx - 1, r) + cell_txy(P, f, 0, r));
    } else {
        if (i == 0) { double a = cell_txy(P, f, 0, r), b = cell_txy(P, f, 1, r); return a - (b - a) * 0.5; }
        if (i == Nx) { double a = cell_txy(P, f, Nx - 1, r), b = cell_txy(P, f, Nx - 2, r); return a + (a - b) * 0.5; }
    }
    return 0.5 * (cell_txy(P, f, i - 1, r) + cell_txy(P, f, i, r));
}
__device__ __forceinline__ double txy_yface(const Params& P, const Cells& f, int c, int j) {
    const int Ny = P.g.Ny;
    if (P.g.py) {
        if (j == 0 || j == Ny) return 0.5 * (cell_txy(P, f, c, Ny - 1) + cell_txy(P, f, c, 0));
    } else {
        if (j == 0) { double a = cell_txy(P, f, c, 0), b = cell_txy(P, f, c, 1); return a - (b - a) * 0.5; }
        if (j == Ny) { double a = cell_txy(P, f, c, Ny - 1), b = cell_txy(P, f, c, Ny - 2); return a + (a - b) * 0.5; }
    }
    return 0.5 * (cell_txy(P, f, c, j - 1) + cell_txy(P, f, c, j));
}

// symmetric_stress_divergence (Operators.jl:620-735) at U face (i,j) and V face (i,j).
__device__ double ssd_x(const Params& P, const Cells& f, int i, int j) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    double dxx;
    if (P.g.px) {
        int ic = (i == Nx) ? 0 : i;
        dxx = (cell_txx(P, f, ic, j) - cell_txx(P, f, wrapi(ic - 1, Nx), j)) * P.g.ihx;
    } else if (i == 0) {
        dxx = (cell_txx(P, f, 1, j) - cell_txx(P, f, 0, j)) * P.g.ihx;
    } else if (i == Nx) {
        dxx = (cell_txx(P, f, Nx - 1, j) - cell_txx(P, f, Nx - 2, j)) * P.g.ihx;
    } else {
        dxx = (cell_txx(P, f, i, j) - cell_txx(P, f, i - 1, j)) * P.g.ihx;
    }
    double dxy;
    if (P.g.py) {
        dxy = (txy_xface(P, f, i, wrapi(j + 1, Ny)) - txy_xface(P, f, i, wrapi(j - 1, Ny))) / (2.0 * P.g.hy);
    } else if (j == 0) {
        dxy = (txy_xface(P, f, i, 1) - txy_xface(P, f, i, 0)) * P.g.ihy;
    } else if (j == Ny - 1) {
        dxy = (txy_xface(P, f, i, Ny - 1) - txy_xface(P, f, i, Ny - 2)) * P.g.ihy;
    } else {
        dxy = (txy_xface(P, f, i, j + 1) - txy_xface(P, f, i, j - 1)) / (2.0 * P.g.hy);
    }
    return dxx + dxy;
}
__device__ double ssd_y(const Params& P, const Cells& f, int i, int j) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    double dyy;
    if (P.g.py) {
        int jc = (j == Ny) ? 0 : j;
        dyy = (cell_tyy(P, f, i, jc) - cell_tyy(P, f, i, wrapi(jc - 1, Ny))) * P.g.ihy;
    } else if (j == 0) {
        dyy = (cell_tyy(P, f, i, 1) - cell_tyy(P, f, i, 0)) * P.g.ihy;
    } else if (j == Ny) {
        dyy = (cell_tyy(P, f, i, Ny - 1) - cell_tyy(P, f, i, Ny - 2)) * P.g.ihy;
    } else {
        dyy = (cell_tyy(P, f, i, j) - cell_tyy(P, f, i, j - 1)) * P.g.ihy;
    }
    double dxy;
    if (P.g.px) {
        dxy = (txy_yface(P, f, wrapi(i + 1, Nx), j) - txy_yface(P, f, wrapi(i - 1, Nx), j)) / (2.0 * P.g.hx);
    } else if (i == 0) {
        dxy = (txy_yface(P, f, 1, j) - txy_yface(P, f, 0, j)) * P.g.ihx;
    } else if (i == Nx - 1) {
        dxy = (txy_yface(P, f, Nx - 1, j) - txy_yface(P, f, Nx - 2, j)) * P.g.ihx;
    } else {
        dxy = (txy_yface(P, f, i + 1, j) - txy_yface(P, f, i - 1, j)) / (2.0 * P.g.hx);
    }
    return dyy + dxy;
}

// Corner velocities for the cross flux u*v (MomentumTransport.jl:60-219).
__device__ __forceinline__ double u_corner(const Params& P, const double* U, int i, int jc) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    int ii = (P.g.px && i == Nx) ? 0 : i;
    if (P.g.py) {
        if (jc == 0 || jc == Ny) return 0.5 * (U[uidx(ii, Ny - 1, Nx)] + U[uidx(ii, 0, Nx)]);
        return 0.5 * (U[uidx(ii, jc - 1, Nx)] + U[uidx(ii, jc, Nx)]);
    }
    if (jc == 0 || jc == Ny) {
        const SideD& s = P.bu.s[jc == 0 ? BOTTOM : TOP];
        if (s.type == EFSI_BC_DIRICHLET) return bval(s, ii);
        double adj = U[uidx(ii, jc == 0 ? 0 : Ny - 1, Nx)];
        return adj + bval(s, ii) * (0.5 * P.g.hy);  // Neumann: linear extension
    }
    return 0.5 * (U[uidx(ii, jc - 1, Nx)] + U[uidx(ii, jc, Nx)]);
}
__device__ __forceinline__ double v_corner(const Params& P, const double* V, int ic, int j) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    int jj = (P.g.py && j == Ny) ? 0 : j;
    if (P.g.px) {
        if (ic == 0 || ic == Nx) return 0.5 * (V[vidx(Nx - 1, jj, Nx)] + V[vidx(0, jj, Nx)]);
        return 0.5 * (V[vidx(ic - 1, jj, Nx)] + V[vidx(ic, jj, Nx)]);
    }
    if (ic == 0 || ic == Nx) {
        const SideD& s = P.bv.s[ic == 0 ? LEFT : RIGHT];
        if (s.type == EFSI_BC_DIRICHLET) return bval(s, jj);
        double adj = V[vidx(ic == 0 ? 0 : Nx - 1, jj, Nx)];
        return adj + bval(s, jj) * (0.5 * P.g.hx);
    }
    return 0.5 * (V[vidx(ic - 1, jj, Nx)] + V[vidx(ic, jj, Nx)]);
}

// Conservative convection minus S*v (MomentumTransport.jl:252-337) at U face (i,j).
__device__ double conv_x(const Params& P, const double* U, const double* V, const double* G, int i, int j) {
    const int Nx = P.g.Nx;
    if (!P.g.px && (i == 0 || i == Nx)) return 0.0;
    int ic = (i == Nx) ? 0 : i;  // periodic duplicate face
    int im = wrapi(ic - 1, Nx);
    auto u2 = [&](int c) {
        double ur = (P.g.px && c == Nx - 1) ? U[uidx(0, j, Nx)] : U[uidx(c + 1, j, Nx)];
        double uc = 0.5 * U[uidx(c, j, Nx)] + 0.5 * ur;
        return uc * uc;
    };
    double cu = (u2(ic) - u2(im)) * P.g.ihx +
                (u_corner(P, U, ic, j + 1) * v_corner(P, V, ic, j + 1) - u_corner(P, U, ic, j) * v_corner(P, V, ic, j)) *
                    P.g.ihy;
    if (G) {
        double Sx = 0.5 * G[cidx(im, j, Nx)] + 0.5 * G[cidx(ic, j, Nx)];
        cu -= Sx * U[uidx(ic, j, Nx)];
    }
    return cu;
}
__device__ double conv_y(const Params& P, const double* U, const double* V, const double* G, int i, int j) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    if (!P.g.py && (j == 0 || j == Ny)) return 0.0;
    int jc = (j == Ny) ? 0 : j;
    int jm = wrapi(jc - 1, Ny);
    auto v2 = [&](int c) {
        double vt = (P.g.py && c == Ny - 1) ? V[vidx(i, 0, Nx)] : V[vidx(i, c + 1, Nx)];
        double vc = 0.5 * V[vidx(i, c, Nx)] + 0.5 * vt;
        return vc * vc;
    };
    double cv = (u_corner(P, U, i + 1, jc) * v_corner(P, V, i + 1, jc) - u_corner(P, U, i, jc) * v_corner(P, V, i, jc)) *
                    P.g.ihx +
                (v2(jc) - v2(jm)) * P.g.ihy;
    if (G) {
        double Sy = 0.5 * G[cidx(i, jm, Nx)] + 0.5 * G[cidx(i, jc, Nx)];
        cv -= Sy * V[vidx(i, jc, Nx)];
    }
    return cv;
}

// scalar_gradient of phi at faces with the phi boundary data (Operators.jl:189-356).
__device__ __forceinline__ double sgrad_x(const Params& P, const BCD& bc, const double* f, int i, int j) {
    const int Nx = P.g.Nx;
    if (P.g.px) {
        int ic = (i == Nx) ? 0 : i;
        return (f[cidx(ic, j, Nx)] - f[cidx(wrapi(ic - 1, Nx), j, Nx)]) * P.g.ihx;
    }
    if (i == 0 || i == Nx) {
        const SideD& s = bc.s[i == 0 ? LEFT : RIGHT];
        double in = f[cidx(i == 0 ? 0 : Nx - 1, j, Nx)];
        double sg = i == 0 ? -1.0 : 1.0, dist = 0.5 * P.g.hx;
        if (bdir(s, j)) return i == 0 ? in / dist - bval(s, j) / dist : bval(s, j) / dist - in / dist;
        if (s.type == EFSI_BC_NEUMANN) return sg * bval(s, j);
        if (s.type == EFSI_BC_MIXED) return sg * bneu(s, j);
        return 0.0;
    }
    return (f[cidx(i, j, Nx)] - f[cidx(i - 1, j, Nx)]) * P.g.ihx;
}
__device__ __forceinline__ double sgrad_y(const Params& P, const BCD& bc, const double* f, int i, int j) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    if (P.g.py) {
        int jc = (j == Ny) ? 0 : j;
        return (f[cidx(i, jc, Nx)] - f[cidx(i, wrapi(jc - 1, Ny), Nx)]) * P.g.ihy;
    }
    if (j == 0 || j == Ny) {
        const SideD& s = bc.s[j == 0 ? BOTTOM : TOP];
        double in = f[cidx(i, j == 0 ? 0 : Ny - 1, Nx)];
        double sg = j == 0 ? -1.0 : 1.0, dist = 0.5 * P.g.hy;
        if (bdir(s, i)) return j == 0 ? in / dist - bval(s, i) / dist : bval(s, i) / dist - in / dist;
        if (s.type == EFSI_BC_NEUMANN) return sg * bval(s, i);
        if (s.type == EFSI_BC_MIXED) return sg * bneu(s, i);
        return 0.0;
    }
    return (f[cidx(i, j, Nx)] - f[cidx(i, j - 1, Nx)]) * P.g.ihy;
}
// interpolate_center_to_{x,y}_faces with constant copy at walls (Operators.jl:110-159).
__device__ __forceinline__ double c2fx(const Params& P, const double* f, int i, int j) {
    const int Nx = P.g.Nx;
    if (i == 0 || i == Nx) {
        if (P.g.px) return 0.5 * f[cidx(Nx - 1, j, Nx)] + 0.5 * f[cidx(0, j, Nx)];
        return f[cidx(i == 0 ? 0 : Nx - 1, j, Nx)];
    }
    return 0.5 * f[cidx(i - 1, j, Nx)] + 0.5 * f[cidx(i, j, Nx)];
}
__device__ __forceinline__ double c2fy(const Params& P, const double* f, int i, int j) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    if (j == 0 || j == Ny) {
        if (P.g.py) return 0.5 * f[cidx(i, Ny - 1, Nx)] + 0.5 * f[cidx(i, 0, Nx)];
        return f[cidx(i, j == 0 ? 0 : Ny - 1, Nx)];
    }
    return 0.5 * f[cidx(i, j - 1, Nx)] + 0.5 * f[cidx(i, j, Nx)];
}

__device__ __forceinline__ double body_x(const Params& P, double t, int j) {  // TransportConstitutive.jl:369-397
    if (P.md.body_force == EFSI_FORCE_CONSTANT) return P.md.body_force_param[0];
    if (P.md.body_force == EFSI_FORCE_KOLMOGOROV) {
        double y = (j + 0.5) * P.g.hy;
        return P.md.body_force_param[0] * sin(P.md.body_force_param[1] * y + P.md.body_force_param[2]);
    }
    return 0.0;
}
__device__ __forceinline__ double body_y(const Params& P) {
    return P.md.body_force == EFSI_FORCE_CONSTANT ? P.md.body_force_param[1] : 0.0;
}

// Interior forms of conv_x/conv_y/ssd_x/ssd_y for 1 <= i <= Nx-2, 1 <= j <= Ny-2: the
// branches the general helpers take at such faces whatever the periodicity, with the
// same arithmetic, so no boundary test is left in the inlined code.
__device__ __forceinline__ double conv_x_in(const Params& P, const double* U, const double* V, const double* G, int i,
                                           int j) {
    const int Nx = P.g.Nx;
    auto u2 = [&](int c) {
        double uc = 0.5 * U[uidx(c, j, Nx)] + 0.5 * U[uidx(c + 1, j, Nx)];
        return uc * uc;
    };
    auto uc = [&](int jc) { return 0.5 * (U[uidx(i, jc - 1, Nx)] + U[uidx(i, jc, Nx)]); };
    auto vc = [&](int jj) { return 0.5 * (V[vidx(i - 1, jj, Nx)] + V[vidx(i, jj, Nx)]); };
    double cu = (u2(i) - u2(i - 1)) * P.g.ihx + (uc(j + 1) * vc(j + 1) - uc(j) * vc(j)) * P.g.ihy;
    if (G) {
        double Sx = 0.5 * G[cidx(i - 1, j, Nx)] + 0.5 * G[cidx(i, j, Nx)];
        cu -= Sx * U[uidx(i, j, Nx)];
    }
    return cu;
}
__device__ __forceinline__ double conv_y_in(const Params& P, const double* U, const double* V, const double* G, int i,
                                           int j) {
    const int Nx = P.g.Nx;
    auto v2 = [&](int c) {
        double vc = 0.5 * V[vidx(i, c, Nx)] + 0.5 * V[vidx(i, c + 1, Nx)];
        return vc * vc;
    };
    auto uc = [&](int ii) { return 0.5 * (U[uidx(ii, j - 1, Nx)] + U[uidx(ii, j, Nx)]); };
    auto vc = [&](int ic) { return 0.5 * (V[vidx(ic - 1, j, Nx)] + V[vidx(ic, j, Nx)]); };
    double cv = (uc(i + 1) * vc(i + 1) - uc(i) * vc(i)) * P.g.ihx + (v2(j) - v2(j - 1)) * P.g.ihy;
    if (G) {
        double Sy = 0.5 * G[cidx(i, j - 1, Nx)] + 0.5 * G[cidx(i, j, Nx)];
        cv -= Sy * V[vidx(i, j, Nx)];
    }
    return cv;
}
__device__ __forceinline__ double ssd_x_in(const Params& P, const Cells& f, int i, int j) {
    auto xface = [&](int r) { return 0.5 * (cell_txy(P, f, i - 1, r) + cell_txy(P, f, i, r)); };
    double dxx = (cell_txx(P, f, i, j) - cell_txx(P, f, i - 1, j)) * P.g.ihx;
    double dxy = (xface(j + 1) - xface(j - 1)) / (2.0 * P.g.hy);
    return dxx + dxy;
}
__device__ __forceinline__ double ssd_y_in(const Params& P, const Cells& f, int i, int j) {
    auto yface = [&](int c) { return 0.5 * (cell_txy(P, f, c, j - 1) + cell_txy(P, f, c, j)); };
    double dyy = (cell_tyy(P, f, i, j) - cell_tyy(P, f, i, j - 1)) * P.g.ihy;
    double dxy = (yface(i + 1) - yface(i - 1)) / (2.0 * P.g.hx);
    return dyy + dxy;
}

// 48 registers at most: five blocks per SM
template <bool FULL>
__global__ void __launch_bounds__(256, 5) k_momentum(Params P, double t, const double* __restrict__ U, const double* __restrict__ V,
                           Cells cells, const double* __restrict__ G, const double* __restrict__ kappa,
                           double* Fx, double* Fy) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const bool elastic = P.md.elastic_stress != EFSI_ELASTIC_NONE ||
                         (P.md.viscosity != EFSI_VISC_NONE && G != nullptr);
    if (i >= 1 && i <= Nx - 2 && j >= 1 && j <= Ny - 2) {
        double fx = -conv_x_in(P, U, V, G, i, j) + body_x(P, t, j);
        double fy = -conv_y_in(P, U, V, G, i, j) + body_y(P);
        if (kappa) {
            fx += P.md.capillary_coefficient * c2fx(P, kappa, i, j) * sgrad_x(P, P.bphi, cells.phi, i, j);
            fy += P.md.capillary_coefficient * c2fy(P, kappa, i, j) * sgrad_y(P, P.bphi, cells.phi, i, j);
        }
        if (elastic) {
            fx += ssd_x_in(P, cells, i, j);
            fy += ssd_y_in(P, cells, i, j);
        }
        Fx[FULL ? uidx(i, j, Nx) : cidx(i, j, Nx)] = fx;
        Fy[FULL ? vidx(i, j, Nx) : cidx(i, j, Nx)] = fy;
        return;
    }
    // x-momentum at U face (i, j)
    if (j < Ny && (FULL ? i <= Nx : i < Nx)) {
        double fx = -conv_x(P, U, V, G, i, j) + body_x(P, t, j);
        if (kappa) fx += P.md.capillary_coefficient * c2fx(P, kappa, i, j) * sgrad_x(P, P.bphi, cells.phi, i, j);
        if (elastic) fx += ssd_x(P, cells, i, j);
        Fx[FULL ? uidx(i, j, Nx) : cidx(i, j, Nx)] = fx;
    }
    if (i < Nx && (FULL ? j <= Ny : j < Ny)) {
        double fy = -conv_y(P, U, V, G, i, j) + body_y(P);
        if (kappa) fy += P.md.capillary_coefficient * c2fy(P, kappa, i, j) * sgrad_y(P, P.bphi, cells.phi, i, j);
        if (elastic) fy += ssd_y(P, cells, i, j);
        Fy[FULL ? vidx(i, j, Nx) : cidx(i, j, Nx)] = fy;
    }
}

void launch_momentum_rhs(const Params& P, double t, const StageFields& f, const double* kappa, double* Eu,
                         double* Ev, DevStatus*, cudaStream_t s) {
    Cells c{f.phi, f.sxx, f.syy, f.sxy, f.G};
    k_momentum<false><<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, t, f.U, f.V, c, f.G, kappa, Eu, Ev);
}
void launch_momentum_full(const Params& P, double t, const StageFields& f, const double* kappa, double* Fx,
                          double* Fy, DevStatus*, cudaStream_t s) {
    Cells c{f.phi, f.sxx, f.syy, f.sxy, f.G};
    k_momentum<true><<<grid2(P.g.Nx + 1, P.g.Ny + 1), dim3(BX, BY), 0, s>>>(P, t, f.U, f.V, c, f.G, kappa, Fx, Fy);
}

// ---- capillarity (Capillarity.jl:96-188): smoothing passes, normals, curvature -------------------
__global__ void k_cap_smooth(Params P, const double* __restrict__ in, double* out) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    if (i >= Nx || j >= Ny) return;
    auto at = [&](int a, int b) {
        a = P.g.px ? wrapi(a, Nx) : min(max(a, 0), Nx - 1);
        b = P.g.py ? wrapi(b, Ny) : min(max(b, 0), Ny - 1);
        return in[cidx(a, b, Nx)];
    };
    out[cidx(i, j, Nx)] = 0.25 * at(i, j) + 0.125 * (at(i + 1, j) + at(i - 1, j) + at(i, j + 1) + at(i, j - 1)) +
                          0.0625 * (at(i + 1, j + 1) + at(i - 1, j + 1) + at(i + 1, j - 1) + at(i - 1, j - 1));
}

// kappa = -div(n) with n interpolated to faces (constant copy at walls).
__device__ __forceinline__ void cap_normal(const Params& P, const double* geo, int i, int j, double& nx, double& ny) {
    double gx = 0.5 * sgrad_x(P, P.bphi, geo, i, j) + 0.5 * sgrad_x(P, P.bphi, geo, i + 1, j);
    double gy = 0.5 * sgrad_y(P, P.bphi, geo, i, j) + 0.5 * sgrad_y(P, P.bphi, geo, i, j + 1);
    double d = sqrt(gx * gx + gy * gy + P.md.capillary_delta_normal * P.md.capillary_delta_normal);
    nx = gx / d;
    ny = gy / d;
}
__global__ void k_cap_curvature(Params P, const double* __restrict__ geo, double* kappa) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    if (i >= Nx || j >= Ny) return;
    auto nxf = [&](int f) {  // x-face f of row j
        int a, b;
        if (f == 0 || f == Nx) {
            if (P.g.px) { a = Nx - 1; b = 0; }
            else { a = b = (f == 0 ? 0 : Nx - 1); }
        } else { a = f - 1; b = f; }
        double n1, m1, n2, m2;
        cap_normal(P, geo, a, j, n1, m1);
        cap_normal(P, geo, b, j, n2, m2);
        return a == b ? n1 : 0.5 * n1 + 0.5 * n2;
    };
    auto nyf = [&](int f) {
        int a, b;
        if (f == 0 || f == Ny) {
            if (P.g.py) { a = Ny - 1; b = 0; }
            else { a = b = (f == 0 ? 0 : Ny - 1); }
        } else { a = f - 1; b = f; }
        double n1, m1, n2, m2;
        cap_normal(P, geo, i, a, n1, m1);
        cap_normal(P, geo, i, b, n2, m2);
        return a == b ? m1 : 0.5 * m1 + 0.5 * m2;
    };
    double div = (nxf(i + 1) - nxf(i)) * P.g.ihx + (nyf(j + 1) - nyf(j)) * P.g.ihy;
    kappa[cidx(i, j, Nx)] = -div;
}

void launch_capillary_curvature(const Params& P, const double* phi, double* smooth_a, double* smooth_b,
                                double* kappa, cudaStream_t s) {
    const double* geo = phi;
    for (int p = 0; p < P.md.capillary_smoothing_passes; ++p) {
        double* out = (p & 1) ? smooth_b : smooth_a;
        k_cap_smooth<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, geo, out);
        geo = out;
    }
    k_cap_curvature<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, geo, kappa);
}

// ---- compact viscous operator application (Operators.jl:929-1083, :1115) ------------------------
// Full MAC arrays seen through the accessor interface of visc_A.
struct MacUV {
    const double* u;
    const double* v;
    int Nx;
    __device__ __forceinline__ double U(int i, int j) const { return u[uidx(i, j, Nx)]; }
    __device__ __forceinline__ double V(int i, int j) const { return v[vidx(i, j, Nx)]; }
};

__global__ void k_viscous_apply(Params P, const double* __restrict__ U, const double* __restrict__ V,
                                const double* __restrict__ phi, double* Iu, double* Iv) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    if (i >= Nx || j >= Ny) return;
    if (i >= 1 && i <= Nx - 2 && j >= 1 && j <= Ny - 2) {
        // interior: no boundary data enters; the same arithmetic as below without its tests
        double au, av;
        if (P.md.viscosity == EFSI_VISC_CONSTANT)
            visc_A<true>(P, MuConst{P.md.viscosity_fluid}, MacUV{U, V, Nx}, i, j, au, av);
        else
            visc_A<true>(P, make_mu(P, phi), MacUV{U, V, Nx}, i, j, au, av);
        Iu[cidx(i, j, Nx)] = au;
        Iv[cidx(i, j, Nx)] = av;
        return;
    }
    MuField mu = make_mu(P, phi);
    const double ihx = P.g.ihx, ihy = P.g.ihy;
    auto u = [&](int a, int b) { return U[uidx(a, b, Nx)]; };
    auto v = [&](int a, int b) { return V[vidx(a, b, Nx)]; };
    auto txx = [&](int c, int r) {
        double nxt = c < Nx - 1 ? u(c + 1, r) : (P.g.px ? u(0, r) : bval(P.bu.s[RIGHT], r));
        return 2.0 * mu.c(c, r) * ((nxt - u(c, r)) * ihx);
    };
    auto tyy = [&](int c, int r) {
        double nxt = r < Ny - 1 ? v(c, r + 1) : (P.g.py ? v(c, 0) : bval(P.bv.s[TOP], c));
        return 2.0 * mu.c(c, r) * ((nxt - v(c, r)) * ihy);
    };
    auto txy = [&](int c, int r) {
        double duy = r > 0 ? (u(c, r) - u(c, r - 1)) * ihy : (P.g.py ? (u(c, 0) - u(c, Ny - 1)) * ihy : 0.0);
        double dvx = c > 0 ? (v(c, r) - v(c - 1, r)) * ihx : (P.g.px ? (v(0, r) - v(Nx - 1, r)) * ihx : 0.0);
        return 2.0 * mu.k(c, r) * (0.5 * duy + 0.5 * dvx);
    };
    double axx = txx(i, j) - (i > 0 ? txx(i - 1, j) : (P.g.px ? txx(Nx - 1, j) : 0.0));
    double axy = -txy(i, j) + (j < Ny - 1 ? txy(i, j + 1) : (P.g.py ? txy(i, 0) : 0.0));
    double au = axx * ihx + axy * ihy;
    double ayx = -txy(i, j) + (i < Nx - 1 ? txy(i + 1, j) : (P.g.px ? txy(0, j) : 0.0));
    double ayy = tyy(i, j) - (j > 0 ? tyy(i, j - 1) : (P.g.py ? tyy(i, Ny - 1) : 0.0));
    double av = ayx * ihx + ayy * ihy;
    if (!P.g.py) {
        if (j == 0 && P.bu.s[BOTTOM].type == EFSI_BC_DIRICHLET) {
            double w = mu.k(i, 0) / (P.g.hy * (0.5 * P.g.hy));
            au += -w * u(i, 0) + w * bval(P.bu.s[BOTTOM], i);
        }
        if (j == Ny - 1 && P.bu.s[TOP].type == EFSI_BC_DIRICHLET) {
            double w = mu.k(i, Ny) / (P.g.hy * (0.5 * P.g.hy));
            au += -w * u(i, Ny - 1) + w * bval(P.bu.s[TOP], i);
        }
    }
    if (!P.g.px) {
        if (i == 0 && P.bv.s[LEFT].type == EFSI_BC_DIRICHLET) {
            double w = mu.k(0, j) / (P.g.hx * (0.5 * P.g.hx));
            av += -w * v(0, j) + w * bval(P.bv.s[LEFT], j);
        }
        if (i == Nx - 1 && P.bv.s[RIGHT].type == EFSI_BC_DIRICHLET) {
            double w = mu.k(Nx, j) / (P.g.hx * (0.5 * P.g.hx));
            av += -w * v(Nx - 1, j) + w * bval(P.bv.s[RIGHT], j);
        }
    }
    Iu[cidx(i, j, Nx)] = au;
    Iv[cidx(i, j, Nx)] = av;
}

void launch_viscous_apply(const Params& P, const double* U, const double* V, const double* phi, double* Iu,
                          double* Iv, cudaStream_t s) {
    k_viscous_apply<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, U, V, phi, Iu, Iv);
}

// ---- upwind conservative advection (InterfaceTransport.jl:83-233, StructureTensor.jl:191-343,
//      ResourceTransport.jl:103-271) ----------------------------------------------------------------
template <bool OUTFLOW>
__device__ __forceinline__ double inflow_state(const SideD& s, int k, double interior, double vel, bool low,
                                               DevStatus* st, int where, int i, int j) {
    if (vel == 0.0) return interior;
    bool inflow = low ? vel > 0.0 : vel < 0.0;
    if (!inflow) return interior;
    if (s.type == EFSI_BC_DIRICHLET) return bval(s, k);
    if (OUTFLOW && s.type == EFSI_BC_ADVECTIVE_OUTFLOW) return bval(s, k);
    raise_err(st, DE_NEUMANN_INFLOW, where, i, j, vel);
    return interior;
}

template <bool OUTFLOW>
__device__ double upwind_rhs(const Params& P, const BCD& bc, const double* U, const double* V, const double* q,
                             int i, int j, DevStatus* st, int where) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    auto fx = [&](int f) {
        if (P.g.px) {
            int fc = (f == Nx) ? 0 : f;
            double u = U[uidx(fc, j, Nx)];
            return u * (u >= 0.0 ? q[cidx(wrapi(fc - 1, Nx), j, Nx)] : q[cidx(fc, j, Nx)]);
        }
        double u = U[uidx(f, j, Nx)];
        if (f == 0) {
            double in = q[cidx(0, j, Nx)];
            double b = inflow_state<OUTFLOW>(bc.s[LEFT], j, in, u, true, st, where, f, j);
            return u * (u >= 0.0 ? b : in);
        }
        if (f == Nx) {
            double in = q[cidx(Nx - 1, j, Nx)];
            double b = inflow_state<OUTFLOW>(bc.s[RIGHT], j, in, u, false, st, where, f, j);
            return u * (u >= 0.0 ? in : b);
        }
        return u * (u >= 0.0 ? q[cidx(f - 1, j, Nx)] : q[cidx(f, j, Nx)]);
    };
    auto fy = [&](int f) {
        if (P.g.py) {
            int fc = (f == Ny) ? 0 : f;
            double v = V[vidx(i, fc, Nx)];
            return v * (v >= 0.0 ? q[cidx(i, wrapi(fc - 1, Ny), Nx)] : q[cidx(i, fc, Nx)]);
        }
        double v = V[vidx(i, f, Nx)];
        if (f == 0) {
            double in = q[cidx(i, 0, Nx)];
            double b = inflow_state<OUTFLOW>(bc.s[BOTTOM], i, in, v, true, st, where, i, f);
            return v * (v >= 0.0 ? b : in);
        }
        if (f == Ny) {
            double in = q[cidx(i, Ny - 1, Nx)];
            double b = inflow_state<OUTFLOW>(bc.s[TOP], i, in, v, false, st, where, i, f);
            return v * (v >= 0.0 ? in : b);
        }
        return v * (v >= 0.0 ? q[cidx(i, f - 1, Nx)] : q[cidx(i, f, Nx)]);
    };
    return -((fx(i + 1) - fx(i)) * P.g.ihx + (fy(j + 1) - fy(j)) * P.g.ihy);
}

// ---- structure tensor (StructureTensor.jl:377-551) ---------------------------------------------
__device__ bool sigma_log_product(double a, double d, double b, double& oxx, double& oyy, double& oxy) {
    double m = 0.5 * (a + d), del = 0.5 * (a - d);
    double r = hypot(del, b);
    double lhi = m + r, llo = m - r;
    if (!(isfinite(llo) && isfinite(lhi) && llo > 0.0)) return false;
    double ghi = lhi * log(lhi), glo = llo * log(llo);
    double scale = fmax(1.0, fabs(m));
    double alpha, beta;
    if (r <= 1.0e-12 * scale) {
        alpha = log(m) + 1.0;
        beta = -m;
    } else {
        double den = lhi - llo;
        alpha = (ghi - glo) / den;
        beta = (lhi * glo - llo * ghi) / den;
    }
    oxx = alpha * a + beta;
    oyy = alpha * d + beta;
    oxy = alpha * b;
    return true;
}

__device__ __forceinline__ double wall_u_at_xc(const SideD& s, int i) { return 0.5 * bval(s, i) + 0.5 * bval(s, i + 1); }

// 64 registers at most: four blocks per SM
__global__ void __launch_bounds__(256, 4) k_structure(Params P, const double* __restrict__ U, const double* __restrict__ V,
                            const double* __restrict__ phi, const double* __restrict__ sxx,
                            const double* __restrict__ syy, const double* __restrict__ sxy,
                            const double* __restrict__ G, double* Exx, double* Eyy, double* Exy, DevStatus* st) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    if (i >= Nx || j >= Ny) return;
    const size_t k = cidx(i, j, Nx);
    const double ihx = P.g.ihx, ihy = P.g.ihy;
    auto Uc = [&](int r) { return 0.5 * U[uidx(i, r, Nx)] + 0.5 * U[uidx(i + 1, r, Nx)]; };
    auto Vc = [&](int c) { return 0.5 * V[vidx(c, j, Nx)] + 0.5 * V[vidx(c, j + 1, Nx)]; };
    double ax, ay, ac, dudy, dvdx;  // Operators.jl:474-583
    if (i >= 1 && i <= Nx - 2 && j >= 1 && j <= Ny - 2) {
        // interior: the branches upwind_rhs and the gradients below take here, whatever
        // the periodicity (same arithmetic), with the face velocities loaded once
        const double ul = U[uidx(i, j, Nx)], ur = U[uidx(i + 1, j, Nx)];
        const double vb = V[vidx(i, j, Nx)], vt = V[vidx(i, j + 1, Nx)];
        auto up = [&](const double* q) {
            auto c = [&](int a, int b) { return q[cidx(a, b, Nx)]; };
            const double fxr = ur * (ur >= 0.0 ? c(i, j) : c(i + 1, j));
            const double fxl = ul * (ul >= 0.0 ? c(i - 1, j) : c(i, j));
            const double fyt = vt * (vt >= 0.0 ? c(i, j) : c(i, j + 1));
            const double fyb = vb * (vb >= 0.0 ? c(i, j - 1) : c(i, j));
            return -((fxr - fxl) * ihx + (fyt - fyb) * ihy);
        };
        ax = up(sxx);
        ay = up(syy);
        ac = up(sxy);
        dudy = (Uc(j + 1) - Uc(j - 1)) / (2.0 * P.g.hy);
        dvdx = (Vc(i + 1) - Vc(i - 1)) / (2.0 * P.g.hx);
    } else {
        ax = upwind_rhs<false>(P, P.bsxx, U, V, sxx, i, j, st, 4);
        ay = upwind_rhs<false>(P, P.bsyy, U, V, syy, i, j, st, 5);
        ac = upwind_rhs<false>(P, P.bsxy, U, V, sxy, i, j, st, 6);
        if (P.g.py) dudy = (Uc(wrapi(j + 1, Ny)) - Uc(wrapi(j - 1, Ny))) / (2.0 * P.g.hy);
        else if (j == 0) {
            const SideD& s = P.bu.s[BOTTOM];
            dudy = s.type == EFSI_BC_DIRICHLET ? (Uc(0) - wall_u_at_xc(s, i)) / (0.5 * P.g.hy) : -wall_u_at_xc(s, i);
        } else if (j == Ny - 1) {
            const SideD& s = P.bu.s[TOP];
            dudy = s.type == EFSI_BC_DIRICHLET ? (wall_u_at_xc(s, i) - Uc(Ny - 1)) / (0.5 * P.g.hy) : wall_u_at_xc(s, i);
        } else dudy = (Uc(j + 1) - Uc(j - 1)) / (2.0 * P.g.hy);
        if (P.g.px) dvdx = (Vc(wrapi(i + 1, Nx)) - Vc(wrapi(i - 1, Nx))) / (2.0 * P.g.hx);
        else if (i == 0) {
            const SideD& s = P.bv.s[LEFT];
            dvdx = s.type == EFSI_BC_DIRICHLET ? (Vc(0) - wall_u_at_xc(s, j)) / (0.5 * P.g.hx) : -wall_u_at_xc(s, j);
        } else if (i == Nx - 1) {
            const SideD& s = P.bv.s[RIGHT];
            dvdx = s.type == EFSI_BC_DIRICHLET ? (wall_u_at_xc(s, j) - Vc(Nx - 1)) / (0.5 * P.g.hx) : wall_u_at_xc(s, j);
        } else dvdx = (Vc(i + 1) - Vc(i - 1)) / (2.0 * P.g.hx);
    }
    const double dudx = (U[uidx(i + 1, j, Nx)] - U[uidx(i, j, Nx)]) * ihx;
    const double dvdy = (V[vidx(i, j + 1, Nx)] - V[vidx(i, j, Nx)]) * ihy;
    const double divv = dudx + dvdy;
    double kxx = 0, kxy = 0, kyx = 0, kyy = 0;
    if (G) growth_K(P.md, G[k], kxx, kxy, kyx, kyy);
    double a11 = dudx - kxx, a12 = dudy - kxy, a21 = dvdx - kyx, a22 = dvdy - kyy;
    double sx = sxx[k], sy = syy[k], sc = sxy[k];
    double dxx = 2.0 * (a11 * sx + a12 * sc);
    double dyy = 2.0 * (a21 * sc + a22 * sy);
    double dxy = a21 * sx + a12 * sy + (a11 + a22) * sc;
    double rxx = 0, ryy = 0, rxy = 0;
    if (P.md.tensor_relaxation == EFSI_RELAX_MAXWELL) {
        double r = P.md.relaxation_rate;
        rxx = -r * (sx - 1.0); ryy = -r * (sy - 1.0); rxy = -r * sc;
    }
    double exx = 0, eyy = 0, exy = 0;
    if (P.nu.structure_extension == EFSI_EXT_GEOMETRIC) {
        double kappa = P.nu.extension_rate * pow(1.0 - clamp01(phi[k]), P.nu.extension_exponent);
        if (kappa != 0.0) {
            double gx, gy, gxy;
            if (sigma_log_product(sx, sy, sc, gx, gy, gxy)) {
                exx = -kappa * gx; eyy = -kappa * gy; exy = -kappa * gxy;
            } else {
                raise_err(st, DE_NON_SPD, 0, i, j, sx);
            }
        }
    }
    Exx[k] = (ax + sx * divv) + dxx + rxx + exx;
    Eyy[k] = (ay + sy * divv) + dyy + ryy + eyy;
    Exy[k] = (ac + sc * divv) + dxy + rxy + exy;
}

void launch_structure_rhs(const Params& P, const StageFields& f, double* Exx, double* Eyy, double* Exy,
                          DevStatus* st, cudaStream_t s) {
    k_structure<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, f.U, f.V, f.phi, f.sxx, f.syy, f.sxy, f.G, Exx,
                                                              Eyy, Exy, st);
}

// ---- resource (ResourceTransport.jl:331-342; Operators.jl:361-384) ---------------------------------
__global__ void k_resource(Params P, const double* __restrict__ U, const double* __restrict__ V,
                           const double* __restrict__ phi, const double* __restrict__ c, double* Ec, double* Ic,
                           DevStatus* st) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    if (i >= Nx || j >= Ny) return;
    const size_t k = cidx(i, j, Nx);
    double sink = 0.0;
    if (P.md.resource_consumption == EFSI_CONSUMPTION_SATURATING) {
        sink = P.md.consumption_rate * phi[k] * c[k] / (P.md.consumption_half_saturation + c[k]);
        if (!isfinite(sink)) raise_err(st, DE_NONFINITE_SINK, 0, i, j, sink);
    }
    Ec[k] = upwind_rhs<true>(P, P.bc, U, V, c, i, j, st, 3) - sink;
    if (Ic) {
        // Div(D_face * scalar_gradient(c)) with D interpolated to faces (copy at walls).
        auto Dc = [&](int a, int b) {
            double d = diffusivity(P.md, phi[cidx(a, b, Nx)]);
            return d;
        };
        auto Dfx = [&](int f) {
            if (f == 0 || f == Nx) {
                if (P.g.px) return 0.5 * Dc(Nx - 1, j) + 0.5 * Dc(0, j);
                return Dc(f == 0 ? 0 : Nx - 1, j);
            }
            return 0.5 * Dc(f - 1, j) + 0.5 * Dc(f, j);
        };
        auto Dfy = [&](int f) {
            if (f == 0 || f == Ny) {
                if (P.g.py) return 0.5 * Dc(i, Ny - 1) + 0.5 * Dc(i, 0);
                return Dc(i, f == 0 ? 0 : Ny - 1);
            }
            return 0.5 * Dc(i, f - 1) + 0.5 * Dc(i, f);
        };
        double dself = Dc(i, j);
        if (!(isfinite(dself) && dself > 0.0)) raise_err(st, DE_BAD_DIFFUSIVITY, 0, i, j, dself);
        Ic[k] = (Dfx(i + 1) * sgrad_x(P, P.bc, c, i + 1, j) - Dfx(i) * sgrad_x(P, P.bc, c, i, j)) * P.g.ihx +
                (Dfy(j + 1) * sgrad_y(P, P.bc, c, i, j + 1) - Dfy(j) * sgrad_y(P, P.bc, c, i, j)) * P.g.ihy;
    }
}

void launch_resource_rhs(const Params& P, const StageFields& f, double* Ec, double* Ic, DevStatus* st,
                         cudaStream_t s) {
    k_resource<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, f.U, f.V, f.phi, f.c, Ec, Ic, st);
}

// ---- final commit and StepReport (TimeIntegrationIMEX.jl:1231-1255) ----------------------------
__global__ void k_finalize(Params P, const double* __restrict__ Us, const double* __restrict__ Vs,
                           const double* __restrict__ phis, const double* __restrict__ cs,
                           const double* __restrict__ sxs, const double* __restrict__ sys,
                           const double* __restrict__ sxys, double* U, double* V, double* phi, double* c, double* sxx,
                           double* syy, double* sxy, double* rep, long long* nonspd, RedSlot rmax, RedSlot rsum,
                           const DevStatus* st) {
    __shared__ double sh[32 * 5];
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const bool ok = st->code == 0;
    if (ok) {
        if (i <= Nx && j < Ny) U[uidx(i, j, Nx)] = Us[uidx(i, j, Nx)];
        if (i < Nx && j <= Ny) V[vidx(i, j, Nx)] = Vs[vidx(i, j, Nx)];
    }
    double mx[5] = {-1e308, -1e308, -1e308, -1e308, -1e308};
    double cnt[1] = {0.0};
    if (i < Nx && j < Ny) {
        size_t k = cidx(i, j, Nx);
        double p = phis[k], r = cs[k], a = sxs[k], d = sys[k], b = sxys[k];
        if (ok) { phi[k] = p; c[k] = r; sxx[k] = a; syy[k] = d; sxy[k] = b; }
        double det = a * d - b * b;
        double lmin = 0.5 * (a + d - hypot(a - d, 2.0 * b));
        mx[0] = -p; mx[1] = p; mx[2] = -r; mx[3] = -lmin; mx[4] = fabs(det - 1.0);
        if (!(isfinite(lmin) && lmin > 0.0)) cnt[0] = 1.0;
    }
    double t5[5], t1[1];
    if (grid_reduce<5, true>(mx, rmax, t5, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        rep[0] = -t5[0]; rep[1] = t5[1]; rep[2] = -t5[2]; rep[3] = -t5[3]; rep[4] = t5[4];
    }
    if (grid_reduce<1, false>(cnt, rsum, t1, sh) && threadIdx.x == 0 && threadIdx.y == 0)
        *nonspd = (long long)llrint(t1[0]);
}

void launch_finalize(const Params& P, const double* Us, const double* Vs, const double* phis, const double* cs,
                     const double* sxs, const double* sys, const double* sxys, double* U, double* V, double* phi,
                     double* c, double* sxx, double* syy, double* sxy, double* report6, long long* nonspd,
                     const RedSlot& rmax, const RedSlot& rsum, const DevStatus* st, cudaStream_t s) {
    k_finalize<<<grid2(P.g.Nx + 1, P.g.Ny + 1), dim3(BX, BY), 0, s>>>(P, Us, Vs, phis, cs, sxs, sys, sxys, U, V, phi,
                                                                     c, sxx, syy, sxy, report6, nonspd, rmax, rsum,
                                                                     st);
}

// ---- |u|_max for dynamic ACDI mobility (PhaseFieldMethods.jl:576-596) -----------------------------
__global__ void k_umax(Params P, const double* __restrict__ U, const double* __restrict__ V, double* out, RedSlot rs) {
    __shared__ double sh[32];
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx;
    double m[1] = {0.0};
    if (i < Nx && j < P.g.Ny) {
        double uc = 0.5 * U[uidx(i, j, Nx)] + 0.5 * U[uidx(i + 1, j, Nx)];
        double vc = 0.5 * V[vidx(i, j, Nx)] + 0.5 * V[vidx(i, j + 1, Nx)];
        m[0] = hypot(uc, vc);
    }
    double t[1];
    if (grid_reduce<1, true>(m, rs, t, sh) && threadIdx.x == 0 && threadIdx.y == 0)
        *out = P.md.pf_param[0] * fmax(t[0], 0.0);
}

void launch_umax(const Params& P, const double* U, const double* V, double* out, const RedSlot& rs,
                 cudaStream_t s) {
    k_umax<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, U, V, out, rs);
}

__global__ void k_copy(double* __restrict__ dst, const double* __restrict__ src, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        dst[k] = src[k];
}
void launch_copy(double* dst, const double* src, size_t n, cudaStream_t s) {
    int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    k_copy<<<blocks, 256, 0, s>>>(dst, src, n);
}

}  // namespace efsi
