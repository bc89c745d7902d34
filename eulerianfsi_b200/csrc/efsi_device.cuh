// efsi_device.cuh — pointwise constitutive closures and the viscosity accessor,
// shared by the explicit kernels and the implicit solvers.
#pragma once

#include "efsi_common.cuh"

namespace efsi {

// ---- constitutive closures (pointwise) ----------------------------------------------------
__device__ __forceinline__ double growth_G(const efsi_models& md, double phi, double c) {  // GrowthModels.jl:214-250
    if (md.growth_source == EFSI_GROWTH_CONSTANT) return md.growth_rate * phi;
    if (md.growth_source == EFSI_GROWTH_SATURATING) return md.growth_rate * phi * c / (md.growth_half_saturation + c);
    return 0.0;
}
__device__ __forceinline__ void growth_K(const efsi_models& md, double G, double& kxx, double& kxy, double& kyx,
                                         double& kyy) {  // GrowthModels.jl:268-318
    if (md.growth_tensor == EFSI_GTENSOR_DIRECTIONAL) {
        double tx = md.growth_direction_x, ty = md.growth_direction_y;
        kxx = tx * tx * G; kxy = tx * ty * G; kyx = tx * ty * G; kyy = ty * ty * G;
    } else {
        kxx = 0.5 * G; kyy = 0.5 * G; kxy = 0.0; kyx = 0.0;
    }
}
__device__ __forceinline__ double viscosity(const efsi_models& md, double phi) {  // TransportConstitutive.jl:131-165
    if (md.viscosity == EFSI_VISC_HARMONIC) {
        double p = clamp01(phi);
        return 1.0 / ((1.0 - p) / md.viscosity_fluid + p / md.viscosity_structure);
    }
    return md.viscosity == EFSI_VISC_CONSTANT ? md.viscosity_fluid : 0.0;
}
__device__ __forceinline__ double diffusivity(const efsi_models& md, double phi) {  // :217-240
    if (md.diffusivity == EFSI_DIFF_HARMONIC)
        return 1.0 / ((1.0 - phi) / md.diffusivity_fluid + phi / md.diffusivity_structure);
    return md.diffusivity == EFSI_DIFF_CONSTANT ? md.diffusivity_fluid : 0.0;
}

// Viscosity accessor: constant, or evaluated from phi (cell centres and the
// bilinear corner values of interpolate_center_to_corners, Operators.jl:162-185).
struct MuField {
    const double* phi;
    int kind;           // EFSI_VISC_*
    double mf, ms;      // fluid / structure viscosity
    int Nx, Ny, px, py;
    __device__ __forceinline__ double c(int i, int j) const {
        if (kind == EFSI_VISC_CONSTANT) return mf;
        if (kind == EFSI_VISC_HARMONIC) {
            double p = clamp01(phi[cidx(i, j, Nx)]);
            return 1.0 / ((1.0 - p) / mf + p / ms);
        }
        return 0.0;
    }
    __device__ double k(int i, int jj) const {
        if (kind == EFSI_VISC_CONSTANT) return mf;
        auto xf = [&](int r) {
            if (px && (i == 0 || i == Nx)) return 0.5 * (c(Nx - 1, r) + c(0, r));
            if (i == 0) return c(0, r);
            if (i == Nx) return c(Nx - 1, r);
            return 0.5 * (c(i - 1, r) + c(i, r));
        };
        if (py && (jj == 0 || jj == Ny)) return 0.5 * (xf(Ny - 1) + xf(0));
        if (jj == 0) return xf(0);
        if (jj == Ny) return xf(Ny - 1);
        return 0.5 * (xf(jj - 1) + xf(jj));
    }
};
__device__ __forceinline__ MuField make_mu(const Params& P, const double* phi) {
    return MuField{phi, P.md.viscosity, P.md.viscosity_fluid, P.md.viscosity_structure, P.g.Nx, P.g.Ny, P.g.px, P.g.py};
}

// Matrix part of the viscous operator (no boundary data), rows u(i,j) and v(i,j).
// INT: (i,j) is at least one cell away from every edge, so no boundary branch is
// taken (the same arithmetic as the general path there, without its tests).
// Constant viscosity known to the compiler (the common case: ConstantViscosity).
struct MuConst {
    double m;
    __device__ __forceinline__ double c(int, int) const { return m; }
    __device__ __forceinline__ double k(int, int) const { return m; }
};

template <bool INT, class X, class MU>
__device__ __forceinline__ void visc_A(const Params& P, const MU& mu, const X& x, int i, int j, double& au,
                                       double& av) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const double ihx = P.g.ihx, ihy = P.g.ihy;
    const bool px = P.g.px, py = P.g.py;
    auto txx = [&](int c, int r) {
        double nxt = (INT || c < Nx - 1) ? x.U(c + 1, r) : (px ? x.U(0, r) : 0.0);
        return 2.0 * mu.c(c, r) * ((nxt - x.U(c, r)) * ihx);
    };
    auto tyy = [&](int c, int r) {
        double nxt = (INT || r < Ny - 1) ? x.V(c, r + 1) : (py ? x.V(c, 0) : 0.0);
        return 2.0 * mu.c(c, r) * ((nxt - x.V(c, r)) * ihy);
    };
    auto txy = [&](int c, int r) {
        double duy = (INT || r > 0) ? (x.U(c, r) - x.U(c, r - 1)) * ihy
                                    : (py ? (x.U(c, 0) - x.U(c, Ny - 1)) * ihy : 0.0);
        double dvx = (INT || c > 0) ? (x.V(c, r) - x.V(c - 1, r)) * ihx
                                    : (px ? (x.V(0, r) - x.V(Nx - 1, r)) * ihx : 0.0);
        return 2.0 * mu.k(c, r) * (0.5 * duy + 0.5 * dvx);
    };
    double axx = txx(i, j) - ((INT || i > 0) ? txx(i - 1, j) : (px ? txx(Nx - 1, j) : 0.0));
    double axy = -txy(i, j) + ((INT || j < Ny - 1) ? txy(i, j + 1) : (py ? txy(i, 0) : 0.0));
    au = axx * ihx + axy * ihy;
    double ayx = -txy(i, j) + ((INT || i < Nx - 1) ? txy(i + 1, j) : (px ? txy(0, j) : 0.0));
    double ayy = tyy(i, j) - ((INT || j > 0) ? tyy(i, j - 1) : (py ? tyy(i, Ny - 1) : 0.0));
    av = ayx * ihx + ayy * ihy;
    if (INT) return;
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

}  // namespace efsi
