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

}  // namespace efsi
